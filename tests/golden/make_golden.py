"""Generate the golden vectors of tests/golden/ by running the reference's own
CUDA code (oracle/_ref, built by `make -C oracle ref` from the reference
sources).  Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py

Cases (seeded synthetic inputs, written with fwi2d_b200.synth):
  A  48 x 96 at 10 m, 20-cell ABC, nt 500, 30 Hz, 3 shots, 24 receivers:
     the harness's seismograms with the source injected in its own launch
     (the golden values), its wavelet, b1d and final fields, and - to record the
     reference's injection race - modeling.exe's and the harness's raw
     forward_solver seismograms;
  B  case A geometry, ABC off, padded velocity = the oracle's random boundary of
     the smoothed model: forward + migration back-propagation
     (inject_seismogram + cross_correlation) and forward + adjoint
     back-propagation (inject_adjoint + build_gradient) of A's seismograms;
  C  37 x 71 at 12.5 m, 13-cell ABC, nt 400, 25 Hz, receivers on row 0:
     modeling.exe seismograms.
Outputs: tests/golden/ref_modeling.npz, ref_backward.npz.
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fwi2d_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = ROOT / "oracle" / "_ref"
OUT = ROOT / "tests" / "golden"


def run(cmd, cwd):
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True, cwd=cwd, timeout=600,
                       env={"TERM": "dumb", "PATH": "/usr/bin:/bin"})
    if r.returncode != 0:
        raise SystemExit(f"{cmd} failed rc={r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r.stdout


def ld(p, n):
    return np.fromfile(p, np.float32, n)


def modeling_case(tmp, tag, **kw):
    """modeling.exe as shipped, then the harness (raw and race-free injection)."""
    case, vp = synth.small_case(Path(tmp) / tag, **kw)
    run([REF / "modeling.exe", case.params], case.root)
    nt, nr = case.nt, len(case.rx)
    us = int(np.float32(1e6) * np.float32(case.dt))
    exe = np.stack([ld(case.root / "data" / f"seismogram_nt{nt}_nr{nr}_{us}us_shot_{s + 1}.bin", nt * nr)
                    .reshape(nr, nt).T for s in range(len(case.sx))])
    h = Path(tmp) / f"h{tag}"
    h.mkdir()
    run([REF / "ref_harness", case.params, h], case.root)
    seis = lambda name: np.stack([ld(h / f"{name}_{s + 1}.bin", nt * nr).reshape(nr, nt).T
                                  for s in range(len(case.sx))])
    return case, vp, exe, seis("seis_raw"), seis("seis"), h


def main():
    if not (REF / "modeling.exe").exists():
        raise SystemExit("oracle/_ref/modeling.exe is missing: run `make -C oracle ref` where the reference is")
    with tempfile.TemporaryDirectory() as tmp:
        # ---- A
        kwA = dict(seed=11)
        caseA, vpA, exeA, rawA, seisA, hA = modeling_case(tmp, "A", **kwA)
        nb = 20
        nzz, nxx = caseA.nz + 2 * nb, caseA.nx + 2 * nb
        wavelet = ld(hA / "wavelet.bin", caseA.nt)
        b1d = ld(hA / "b1d.bin", nb)
        p1 = ld(hA / "p_1.bin", nzz * nxx).reshape(nxx, nzz).T
        pold1 = ld(hA / "pold_1.bin", nzz * nxx).reshape(nxx, nzz).T
        # ---- C
        kwC = dict(seed=13, nz=37, nx=71, dh=12.5, nt=400, fmax=25.0, nshots=2, nrec=15, boundary=150.0)
        caseC, vpC, exeC, rawC, seisC, _ = modeling_case(tmp, "C", **kwC)
        np.savez_compressed(OUT / "ref_modeling.npz", A_kwargs=repr(kwA), A_seis=seisA, A_seis_exe=exeA,
                            A_seis_raw=rawA, A_wavelet=wavelet, A_b1d=b1d, A_p1=p1, A_pold1=pold1,
                            C_kwargs=repr(kwC), C_seis=seisC, C_seis_exe=exeC)
        # ---- B
        smooth = synth.smooth_model(vpA, caseA.dh, 40.0)
        base = O.expand(smooth, nb)
        seed, varVp, ratio = 3, 500.0, 60.0
        bt = O.bumps(nxx, nzz, nb, caseA.dh, ratio, varVp, seed, 0)
        vel = O.rbc(base, nb, caseA.dh, varVp, float(smooth.min()), float(smooth.max()), seed, 0, bt)
        np.ascontiguousarray(vel.T).tofile(Path(tmp) / "vel.bin")
        for s in range(len(caseA.sx)):
            np.ascontiguousarray(seisA[s].T).tofile(Path(tmp) / f"data_{s + 1}.bin")
        hB = Path(tmp) / "hB"
        hB.mkdir()
        run([REF / "ref_harness", caseA.params, hB, Path(tmp) / "vel.bin", str(Path(tmp) / "data_")], caseA.root)
        acc = {}
        for tag in ("image", "image_illum", "grad", "grad_illum"):
            acc[tag] = np.stack([ld(hB / f"{tag}_{s + 1}.bin", nzz * nxx).reshape(nxx, nzz).T
                                 for s in range(len(caseA.sx))])
        seisB = np.stack([ld(hB / f"seis_{s + 1}.bin", caseA.nt * len(caseA.rx)).reshape(len(caseA.rx), caseA.nt).T
                          for s in range(len(caseA.sx))])
        np.savez_compressed(OUT / "ref_backward.npz", kwargs=repr(kwA), vel=vel, seis_rbc=seisB,
                            **{k: v for k, v in acc.items()})
    print("golden vectors written to", OUT)


if __name__ == "__main__":
    main()
