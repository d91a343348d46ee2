"""The random boundary's draws against the reference's own sampler (CPU).

The reference's random boundary (set_random_boundary, modeling.cu:431-465) is
unseeded, so it cannot be matched draw for draw.  This project keeps its
structure with a seeded counter-based generator (the oracle and the engine are
bit-identical, tests/test_host.py and the GPU tests).  Here that generator is
held to the reference at the level of distributions:

* Poisson-disk point sets: the counts before and after the band filter and the
  nearest-neighbour distances of 64 seeds of the project's sampler against 64
  runs of the reference's poissonDiskSampling (admin.cpp:115-206, run
  unchanged with its std::mt19937 reseeded; tests/golden/ref_pds_stats.json,
  made by tests/golden/make_pds_stats.py), on three geometries;
* bump parameters against the ranges modeling.cu:458-461 draws from:
  r ~ U(0.2 ratio, ratio), A ~ U(0.5 varVp, varVp), sign + with
  probability 1/3 (rand() % 3 == 0).
"""
import json
import math
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from make_pds_stats import GEOMETRIES, point_stats  # noqa: E402

REF = json.loads((GOLDEN / "ref_pds_stats.json").read_text())


@pytest.fixture(scope="module", params=[g[0] for g in GEOMETRIES])
def both(request):
    name, nxx, nzz, dh, nb, ratio = next(g for g in GEOMETRIES if g[0] == request.param)
    x_max, z_max = np.float32((nxx - 1) * dh), np.float32((nzz - 1) * dh)
    ours = [point_stats(O.pds(float(x_max), float(z_max), ratio, seed, 0), float(x_max), float(z_max), nb * dh)
            for seed in range(64)]
    return name, REF["geometries"][name]["per_seed"], ours, ratio


@pytest.mark.parametrize("key", ["n", "kept", "nn_min", "nn_mean", "nn_p90"])
def test_point_set_statistics_match_reference_sampler(both, key):
    """Means over 64 seeds agree within 4 standard errors of their difference."""
    name, ref, ours, _ = both
    a = np.array([r[key] for r in ref], np.float64)
    b = np.array([r[key] for r in ours], np.float64)
    se = math.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    assert abs(a.mean() - b.mean()) <= 4.0 * se, (name, key, a.mean(), b.mean(), se)


def test_spread_of_point_counts_matches(both):
    """The seed-to-seed spread of the point count agrees within a factor 1.6."""
    name, ref, ours, _ = both
    sa = np.std([r["n"] for r in ref], ddof=1)
    sb = np.std([r["n"] for r in ours], ddof=1)
    assert 1 / 1.6 < sb / sa < 1.6, (name, sa, sb)


def test_bump_parameter_ranges_and_sign_ratio():
    ratio, var = 200.0, 500.0
    t = np.concatenate([O.bumps(701, 351, 100, 10.0, ratio, var, seed, s) for seed in range(4) for s in range(4)])
    r, A, sign = t[:, 2], t[:, 3], t[:, 4]
    n = len(t)
    assert n > 2000
    assert r.min() >= 0.2 * ratio and r.max() < ratio
    assert A.min() >= 0.5 * var and A.max() < var
    # uniform: mean at the middle of the range within 4 standard errors
    assert abs(r.mean() - 0.6 * ratio) < 4 * (0.8 * ratio / math.sqrt(12 * n))
    assert abs(A.mean() - 0.75 * var) < 4 * (0.5 * var / math.sqrt(12 * n))
    assert set(np.unique(sign)) == {-1.0, 1.0}
    p = float((sign > 0).mean())
    assert abs(p - 1 / 3) < 4 * math.sqrt((1 / 3) * (2 / 3) / n), p
