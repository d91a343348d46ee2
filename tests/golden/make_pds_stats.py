"""Statistics of the reference's own Poisson-disk sampler for tests/golden/.

The reference places the Gaussian bumps of its random boundary at the points of
poissonDiskSampling (src/admin/admin.cpp:115-206) that lie outside the inner
box shrunk by half the boundary width (src/modeling/modeling.cu:438-448).  It
draws from an unseeded global std::mt19937, so no run of it can be reproduced;
oracle/_ref/ref_pds (oracle/ref_pds.cpp, built by `make -C oracle ref REF=...`
from the reference sources) reseeds that generator and runs the sampler
unchanged.  This script runs it for 64 seeds on three geometries and records,
per seed, the number of points, the number kept by the band filter and
nearest-neighbour distances, so tests/test_rbc_stats.py can hold this
project's counter-based sampler to the reference's point-set statistics
without the reference present.  Runs on the CPU, from the repository root:

    python tests/golden/make_pds_stats.py
Output: tests/golden/ref_pds_stats.json
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
EXE = ROOT / "oracle" / "_ref" / "ref_pds"
OUT = ROOT / "tests" / "golden" / "ref_pds_stats.json"

# (name, nxx, nzz, dh, nb, ratio): the random boundaries of the benchmark RTM
# geometry, of the FWI survey and of the small parity case
GEOMETRIES = [("rtm_351x701", 701, 351, 10.0, 100, 200.0), ("fwi_501x1901", 1901, 501, 10.0, 100, 200.0),
              ("small_88x136", 136, 88, 10.0, 20, 60.0)]
SEEDS = range(1, 65)


def point_stats(pts: np.ndarray, x_max: float, z_max: float, fnb: float) -> dict:
    """Counts and nearest-neighbour distances of one point set (n, 2)."""
    x, z = pts[:, 0].astype(np.float64), pts[:, 1].astype(np.float64)
    inner = (pts[:, 0] > np.float32(0.5) * np.float32(fnb)) & (pts[:, 0] < np.float32(x_max) - np.float32(0.5) * np.float32(fnb)) & \
            (pts[:, 1] > np.float32(0.5) * np.float32(fnb)) & (pts[:, 1] < np.float32(z_max) - np.float32(0.5) * np.float32(fnb))
    d = np.hypot(x[:, None] - x[None, :], z[:, None] - z[None, :])
    np.fill_diagonal(d, np.inf)
    nn = d.min(1)
    return {"n": int(len(pts)), "kept": int((~inner).sum()), "nn_min": float(nn.min()), "nn_mean": float(nn.mean()),
            "nn_p90": float(np.percentile(nn, 90))}


def main() -> None:
    if not EXE.exists():
        raise SystemExit("oracle/_ref/ref_pds is missing: run `make -C oracle ref REF=<reference checkout>`")
    res = {"source": "oracle/_ref/ref_pds: src/admin/admin.cpp poissonDiskSampling, std::mt19937 reseeded per run",
           "geometries": {}}
    for name, nxx, nzz, dh, nb, ratio in GEOMETRIES:
        x_max, z_max = np.float32((nxx - 1) * dh), np.float32((nzz - 1) * dh)
        rows = []
        for seed in SEEDS:
            r = subprocess.run([str(EXE), str(seed), repr(float(x_max)), repr(float(z_max)), repr(ratio)],
                               capture_output=True, text=True, check=True)
            pts = np.array([[float(v) for v in ln.split()] for ln in r.stdout.splitlines()], np.float32)
            rows.append(point_stats(pts, float(x_max), float(z_max), nb * dh))
        res["geometries"][name] = {"nxx": nxx, "nzz": nzz, "dh": dh, "nb": nb, "ratio": ratio,
                                   "seeds": list(SEEDS), "per_seed": rows}
        n = np.array([r["n"] for r in rows])
        print(f"{name}: points {n.mean():.1f} +- {n.std():.1f}, kept {np.mean([r['kept'] for r in rows]):.1f}")
    OUT.write_text(json.dumps(res, indent=1) + "\n")


if __name__ == "__main__":
    sys.exit(main())
