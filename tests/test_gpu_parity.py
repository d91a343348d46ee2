"""CUDA path vs the CPU oracle on small seeded surveys (run on a B200: -m gpu).

Tolerances: the engine computes in FP32; its outputs are compared with the FP64
oracle (orc_*, liboracle64) and with the oracle's restatement of the
reference's own float arithmetic (liboracle32).  The bar is relative L2 error
below 1e-4 (RTOL); indices and the random-boundary field are bit-exact.
"""
import os
import subprocess

import numpy as np
import pytest

from fwi2d_b200 import api, synth
from fwi2d_b200 import build as B
from oracle import oracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu
RTOL = 1e-4


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    c, vp = synth.small_case(tmp_path_factory.mktemp("small"))
    return c, vp


def _oracle_setup(c, nb):
    wav, tlag = O.wavelet(c.nt, c.dt, c.fmax)
    sx = O.indices(c.sx, c.dh, nb)
    sz = O.indices(c.sz, c.dh, nb)
    rx = O.indices(c.rx, c.dh, nb)
    rz = O.indices(c.rz, c.dh, nb)
    return wav, tlag, sx, sz, rx, rz


def _oracle_modeling(c, vp, nb, factor, bits=64):
    wav, tlag, sx, sz, rx, rz = _oracle_setup(c, nb)
    vel = O.expand(vp, nb)
    tab = O.b1d(nb, factor)
    return [O.forward(vel, nb, tab, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz, bits=bits)[0]
            for s in range(len(c.sx))]


# ---------------------------------------------------------------------------------- modeling
def test_indices_and_wavelet(case):
    c, vp = case
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        d = ctx.dims
        assert d.nb == 20 and d.nzz == c.nz + 40 and d.nxx == c.nx + 40 and d.ldz % 32 == 0
        for s in range(len(c.sx)):
            sx, sz, rx, rz = ctx.indices(s)
            assert sx == O.indices(c.sx[s:s + 1], c.dh, 20)[0] and sz == O.indices(c.sz[s:s + 1], c.dh, 20)[0]
            assert np.array_equal(rx, O.indices(c.rx, c.dh, 20)) and np.array_equal(rz, O.indices(c.rz, c.dh, 20))
        w = ctx.wavelet()
        assert np.array_equal(w, api.util_wavelet(c.nt, c.dt, c.fmax)[0])


def test_modeling_survey_vs_oracle(case):
    c, vp = case
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        seis = ctx.model_survey()
    ref64 = _oracle_modeling(c, vp, 20, 0.004, 64)
    ref32 = _oracle_modeling(c, vp, 20, 0.004, 32)
    for s in range(len(c.sx)):
        e64 = rel_l2(seis[s], ref64[s])
        e32 = rel_l2(seis[s], ref32[s])
        assert e64 < RTOL, (s, e64)
        assert e32 < RTOL, (s, e32)
        assert np.all(seis[s][0] == 0.0)  # sample 0 is never recorded (modeling.cu:347-353)


def test_single_shot_equals_batched_survey(case):
    c, _ = case
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        allv = ctx.model_survey()
        one = ctx.model_shot(1)
    assert np.array_equal(one, allv[1])


def test_set_model_and_cfl(case):
    c, vp = case
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        ctx.set_model(vp * 1.01)
        assert np.array_equal(ctx.get_model(), (vp * 1.01).astype(np.float32))
        with pytest.raises(api.FwiError) as e:
            ctx.set_model(np.full_like(vp, 9000.0))
        assert e.value.code == -4
        with pytest.raises(api.FwiError) as e:
            bad = vp.copy()
            bad[3, 4] = np.nan
            ctx.set_model(bad)
        assert e.value.code == -1


VARIANTS = ["simple", "tma:1,32,2", "tma:1,32,3", "tma:1,16,3", "tma:1,16,4", "tma:2,32,2", "tma:2,16,2",
            "tma:2,16,3", "loop:32,2", "loop:16,3", "loop:16,2", "loop:16,2,3", "resident"]


@pytest.mark.parametrize("nt", [500, 501])  # nt + tlag odd (T = 2 ends with a one-level launch) and even
@pytest.mark.parametrize("variant", VARIANTS)
def test_forward_kernel_variants_vs_oracle(tmp_path, variant, nt):
    c, vp = synth.small_case(tmp_path, nt=nt, fwd_kernel=variant)
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        seis = ctx.model_survey()
    ref = _oracle_modeling(c, vp, 20, 0.004, 64)
    for s in range(len(c.sx)):
        assert rel_l2(seis[s], ref[s]) < RTOL, (variant, s)
        assert np.all(seis[s][0] == 0.0)


def test_forward_variants_agree_on_wide_grid(tmp_path):
    """Several tiles per column and per shot, receivers across tile borders."""
    outs = {}
    for v in ("simple", "tma:1,32,2", "tma:2,16,2", "tma:2,32,2", "loop:32,2", "loop:16,3", "loop:16,2,3", "resident"):
        c, vp = synth.small_case(tmp_path / v.replace(":", "_").replace(",", "_"), nz=260, nx=300, nt=300,
                                 nshots=4, nrec=77, fwd_kernel=v)
        with api.Context(c.params, api.MODE_MODELING) as ctx:
            outs[v] = ctx.model_survey()
    base = outs["simple"]
    for v, o in outs.items():
        assert rel_l2(o, base) < 1e-5, v


def test_resident_kernel_on_benchmark_survey(tmp_path):
    """The benchmark survey's geometry (11 shots of 351 x 701 with the ABC):
    the resident kernel splits every shot over 13 CTAs that exchange halos
    every level; it must agree with the streaming multi-level kernel."""
    outs = {}
    for v in ("loop:16,3", "resident"):
        c, _ = synth.modeling_survey(tmp_path / v.replace(":", "_").replace(",", "_"), seed=0, nt=400, fwd_kernel=v)
        with api.Context(c.params, api.MODE_MODELING) as ctx:
            outs[v] = ctx.model_survey()
            assert ctx.describe().startswith(v.split(":")[0]), ctx.describe()
    assert rel_l2(outs["resident"], outs["loop:16,3"]) < 1e-5


def test_resident_kernel_migration_on_benchmark_geometry(tmp_path):
    """RTM of the benchmark geometry: the forward through the random boundary
    runs with a velocity per shot; the resident and the streaming forward
    kernels (same backward kernel) must give the same image."""
    imgs = {}
    data = None
    for v in ("loop:16,3", "resident"):
        c, vp = synth.modeling_survey(tmp_path / v.replace(":", "_").replace(",", "_"), seed=0, nt=300, fwd_kernel=v,
                              bwd_kernel="loop:16,3")
        if data is None:
            with api.Context(c.params, api.MODE_MODELING) as ctx:
                data = ctx.model_survey()
        with api.Context(c.params, api.MODE_MIGRATION) as ctx:
            ctx.set_model(synth.smooth_model(vp, c.dh, 150.0))
            ctx.rtm_reset()
            ctx.rtm_survey(data)
            imgs[v] = ctx.rtm_raw()[0]
            assert ctx.describe().startswith(v.split(":")[0]), ctx.describe()
    assert rel_l2(imgs["resident"], imgs["loop:16,3"]) < 1e-5


def test_resident_kernel_refuses_a_survey_that_does_not_fit(tmp_path):
    """A column of more than 384 padded rows does not fit the resident kernel's
    tables: asked for it explicitly, the context fails with FWI_ERR_PARAM."""
    c, _ = synth.small_case(tmp_path, nz=380, nx=64, nt=50, nshots=1, nrec=8, fwd_kernel="resident")
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        with pytest.raises(api.FwiError) as e:
            ctx.model_survey()
    assert e.value.code == -1


# ---------------------------------------------------------------------------- random boundary
def test_random_boundary_bit_exact(case):
    c, vp = case
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        d = ctx.dims
        nb = d.rbc_nb
        base = O.expand(vp, nb)
        for seed in (0, 99):
            ctx.set_seed(seed)
            for s in range(len(c.sx)):
                gpu = ctx.random_boundary(s)
                bt = O.bumps(base.shape[1], base.shape[0], nb, c.dh, 60.0, 500.0, seed, s)
                ref = O.rbc(base, nb, c.dh, 500.0, float(vp.min()), float(vp.max()), seed, s, bt)
                assert np.array_equal(gpu, ref), (seed, s, np.abs(gpu - ref).max())


# ------------------------------------------------------------------------------------ migration
def _rtm_data(c, vp):
    return np.stack(_oracle_modeling(c, vp, 20, 0.004, 64)).astype(np.float32)


@pytest.mark.parametrize("variant,bwd", [("auto", "auto"), ("simple", "simple"), ("tma:2,16,2", "loop:16,3"),
                                         ("tma:1,32,2", "loop:16,2"), ("loop:16,2", "loop:8,4"),
                                         ("loop:32,2", "loop:8,3"), ("resident", "loop:8,3")])
def test_rtm_vs_oracle(case, tmp_path, variant, bwd):
    c0, vp = case
    c, _ = synth.small_case(tmp_path, fwd_kernel=variant, bwd_kernel=bwd)
    smooth = synth.smooth_model(vp, c.dh, 40.0)
    data = _rtm_data(c, vp)
    with api.Context(c.params, api.MODE_MIGRATION) as ctx:
        ctx.set_model(smooth)
        nb = ctx.dims.rbc_nb
        vels = [ctx.random_boundary(s) for s in range(len(c.sx))]
        ctx.rtm_reset()
        ctx.rtm_survey(data)
        img, ill = ctx.rtm_raw()
        image = ctx.rtm_image()
    wav, tlag, sx, sz, rx, rz = _oracle_setup(c, nb)
    acc = np.zeros_like(vels[0], np.float64)
    illum = np.zeros_like(acc)
    for s in range(len(c.sx)):
        _, P, Po = O.forward(vels[s], nb, None, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz, bits=64)
        a, b = O.backward(vels[s], data[s], c.nt, tlag, c.dt, c.dh, rx, rz, P, Po, gradient=False, bits=64)
        acc += a
        illum += b
    ref_img, ref_ill = O.crop(acc, nb), O.crop(illum, nb)
    assert rel_l2(img, ref_img) < RTOL
    assert rel_l2(ill, ref_ill) < RTOL
    # Migration::export_seismic (migration.cu:90-115): the post-processing of the
    # engine's own raw image (FP32, as the reference), and the whole section
    # against the FP64 post-processing of the FP64 oracle's raw image.
    idh2 = 1.0 / c.dh**2
    assert rel_l2(image, O.image_post(img, ill, idh2)) < 1e-6
    q = ref_img / ref_ill
    post64 = np.zeros_like(q)
    post64[1:-1] = -(q[:-2] - 2.0 * q[1:-1] + q[2:]) * idh2
    assert rel_l2(image, post64) < RTOL


# ------------------------------------------------------------------------------------ inversion
@pytest.fixture(scope="module")
def fwi_state(case):
    c, vp = case
    init = synth.smooth_model(vp, c.dh, 40.0)
    obs = _rtm_data(c, vp)
    ctx = api.Context(c.params, api.MODE_INVERSION)
    ctx.set_model(init)
    ctx.set_observed(obs)
    nb = ctx.dims.rbc_nb
    vels = [ctx.random_boundary(s) for s in range(len(c.sx))]
    sum_res = ctx.compute_gradient(True)
    graw, gill = ctx.gradient_raw()
    g = ctx.gradient()
    yield dict(c=c, vp=vp, init=init, obs=obs, ctx=ctx, nb=nb, vels=vels, sum_res=sum_res, graw=graw, gill=gill, g=g)
    ctx.close()


def test_misfit_and_gradient_vs_oracle(fwi_state):
    st = fwi_state
    c, init, obs, nb = st["c"], st["init"], st["obs"], st["nb"]
    cal = _oracle_modeling(c, init, 20, 0.004, 64)
    res = [obs[s].astype(np.float64) - cal[s] for s in range(len(c.sx))]
    ref_sum = sum(float((r * r).sum()) for r in res)
    assert abs(st["sum_res"] - ref_sum) / ref_sum < RTOL
    wav, tlag, sx, sz, rx, rz = _oracle_setup(c, nb)
    acc = np.zeros_like(st["vels"][0], np.float64)
    ill = np.zeros_like(acc)
    for s in range(len(c.sx)):
        _, P, Po = O.forward(st["vels"][s], nb, None, wav, c.nt, tlag, c.dt, c.dh, (sx[s], sz[s]), rx, rz, bits=64)
        a, b = O.backward(st["vels"][s], res[s].astype(np.float32), c.nt, tlag, c.dt, c.dh, rx, rz, P, Po,
                          gradient=True, bits=64)
        acc += a
        ill += b
    ref_g, ref_ill = O.crop(acc, nb), O.crop(ill, nb)
    assert rel_l2(st["graw"], ref_g) < RTOL
    assert rel_l2(st["gill"], ref_ill) < RTOL
    post = O.gradient_post(st["graw"], st["gill"], 1.0 / c.dh**2, int(float(c.keys["depth_mask"]) / c.dh))
    assert rel_l2(st["g"], post) < 1e-5
    assert abs(np.abs(st["g"]).max() - 1.0) < 1e-6


@pytest.mark.parametrize("bwd", ["simple", "loop:16,3", "loop:16,2", "loop:8,4", "loop:8,3"])
def test_gradient_backward_variants_agree(fwi_state, tmp_path, bwd):
    """Every backward kernel gives the raw gradient of the fixture (auto plan)."""
    st = fwi_state
    c, _ = synth.small_case(tmp_path, bwd_kernel=bwd)
    with api.Context(c.params, api.MODE_INVERSION) as ctx:
        ctx.set_model(st["init"])
        ctx.set_observed(st["obs"])
        assert abs(ctx.compute_gradient(True) - st["sum_res"]) <= 1e-12 * st["sum_res"]
        g, ill = ctx.gradient_raw()
    assert rel_l2(g, st["graw"]) < 1e-5, bwd
    assert rel_l2(ill, st["gill"]) < 1e-5, bwd


def test_linesearch_optimization_update(fwi_state):
    st = fwi_state
    c, ctx, init = st["c"], st["ctx"], st["init"]
    g = st["g"].astype(np.float32)
    m = (1.0 / (init.astype(np.float32) * init.astype(np.float32))).astype(np.float32)
    d = ctx.dims
    alpha = np.float32(0.02) * (np.float32(1) / (np.float32(d.vmin) ** 2) - np.float32(1) / (np.float32(d.vmax) ** 2))
    f1 = ctx.linesearch_trial(float(alpha))
    trial = (np.float32(1.0) / np.sqrt(m - alpha * g)).astype(np.float32)
    cal = _oracle_modeling(c, trial, 20, 0.004, 64)
    ref = sum(float(((st["obs"][s] - cal[s]) ** 2).sum()) for s in range(len(c.sx)))
    assert abs(f1 - ref) / ref < RTOL
    f0 = float(np.sqrt(np.float32(st["sum_res"])))
    step = ctx.optimization(f0)
    assert np.isfinite(step)
    vnew = ctx.update_model(step)
    mref = m - np.float32(step) * g
    assert rel_l2(vnew, 1.0 / np.sqrt(mref)) < 1e-6
    assert np.array_equal(ctx.get_model(), vnew)


# ---------------------------------------------------------------------------------- executables
def test_modeling_executable_writes_reference_files(case):
    c, vp = case
    r = subprocess.run([str(B.BIN / "modeling"), str(c.params)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Run time:" in r.stdout
    with api.Context(c.params, api.MODE_MODELING) as ctx:
        seis = ctx.model_survey()
    for s in range(len(c.sx)):
        f = c.root / "data" / f"seismogram_nt{c.nt}_nr{len(c.rx)}_1000us_shot_{s + 1}.bin"
        arr = np.fromfile(f, np.float32).reshape(len(c.rx), c.nt).T
        assert np.array_equal(arr, seis[s])


def test_migration_and_inversion_executables(case, tmp_path):
    c, vp = case
    data = _rtm_data(c, vp)
    for s in range(len(c.sx)):
        np.ascontiguousarray(data[s].T).tofile(c.root / "data" / f"input_RTM_{s + 1}.bin")
        np.ascontiguousarray(data[s].T).tofile(
            c.root / "data" / f"seismogram_nt{c.nt}_nr{len(c.rx)}_1000us_shot_{s + 1}.bin")
    init = synth.smooth_model(vp, c.dh, 40.0)
    np.ascontiguousarray(init.T).tofile(c.root / "model.bin")
    r = subprocess.run([str(B.BIN / "migration"), str(c.params)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    img = np.fromfile(c.root / "out" / f"RTM_section_30Hz_{c.nz}x{c.nx}_10m.bin", np.float32)
    assert img.size == c.nz * c.nx and np.isfinite(img).all() and np.abs(img).max() > 0
    r = subprocess.run([str(B.BIN / "inversion"), str(c.params)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    conv = np.loadtxt(c.root / "out" / "convergence_2_iterations.txt")
    assert conv.shape == (3,) and conv[-1] < conv[0]
    for it in (1, 2):
        m = np.fromfile(c.root / "out" / f"model_FWI_iteration_{it}_30Hz_{c.nz}x{c.nx}_10m.bin", np.float32)
        assert m.size == c.nz * c.nx and np.isfinite(m).all()
    fin = np.fromfile(c.root / "out" / f"final_model_FWI_30Hz_{c.nz}x{c.nx}_10m.bin", np.float32)
    assert np.array_equal(fin, np.fromfile(c.root / "out" / f"model_FWI_iteration_2_30Hz_{c.nz}x{c.nx}_10m.bin",
                                           np.float32))


def test_graphs_and_direct_launches_agree(case):
    c, _ = case
    code = ("import sys, numpy as np; sys.path.insert(0, '.'); from fwi2d_b200 import api; "
            f"ctx = api.Context('{c.params}', 0); np.save(sys.argv[1], ctx.model_survey())")
    outs = []
    for env_extra, name in (({}, "a.npy"), ({"FWI2D_NO_GRAPHS": "1"}, "b.npy")):
        env = dict(os.environ, **env_extra)
        p = c.root / name
        r = subprocess.run(["python", "-c", code, str(p)], env=env, capture_output=True, text=True, timeout=300,
                           cwd=str(B.ROOT))
        assert r.returncode == 0, r.stderr
        outs.append(np.load(p))
    assert np.array_equal(outs[0], outs[1])
