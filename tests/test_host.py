"""Host-side set-up of the engine against the reference's rules and the oracle (CPU only)."""
import numpy as np
import pytest
from scipy.special import ndtri

from fwi2d_b200 import api
from oracle import oracle as O


# ---- parameters.txt (admin.cpp:53-98) -------------------------------------------------------
def _pfile(tmp_path, text):
    p = tmp_path / "p.txt"
    p.write_text(text)
    return p


def test_parameter_first_prefix_match_wins(tmp_path):
    p = _pfile(tmp_path, "# x_samples = 1\n x_samples = 2\nx_samples = 201     \nx_samples = 7\n")
    assert api.util_parameter(p, "x_samples") == "201"


def test_parameter_prefix_semantics(tmp_path):
    # the reference matches the key as a prefix of the line (find(target) == 0)
    p = _pfile(tmp_path, "abc_length_extra = 5\nabc_length = 1250\n")
    assert api.util_parameter(p, "abc_length") == "5"


def test_parameter_comment_and_spaces_stripped(tmp_path):
    p = _pfile(tmp_path, "model_file = ../inputs/models/a b.bin   # comment\n")
    assert api.util_parameter(p, "model_file") == "../inputs/models/ab.bin"


def test_parameter_value_starts_two_after_equals(tmp_path):
    p = _pfile(tmp_path, "dt =1e-3\n")
    assert api.util_parameter(p, "dt") == "e-3"


def test_parameter_missing_key_is_param_error(tmp_path):
    p = _pfile(tmp_path, "x = 1\n")
    with pytest.raises(api.FwiError) as e:
        api.util_parameter(p, "z_samples")
    assert e.value.code == -1


def test_parameter_missing_file_is_io_error(tmp_path):
    with pytest.raises(api.FwiError) as e:
        api.util_parameter(tmp_path / "none.txt", "x")
    assert e.value.code == -2


def test_parameter_quote_squeeze_keeps_tail(tmp_path):
    # std::remove without erase (admin.cpp:65-73): kept chars shift left, the tail stays
    p = _pfile(tmp_path, 'name = "ab"\n')
    assert api.util_parameter(p, "name") == 'abb"'


# ---- wavelet (modeling.cu:32-90) -------------------------------------------------------------
@pytest.mark.parametrize("nt,dt,fmax,tlag", [(3001, 1e-3, 30.0, 119), (4001, 1e-3, 15.0, 237), (2001, 1e-3, 50.0, 71)])
def test_wavelet_tlag_and_filter(nt, dt, fmax, tlag):
    w, tl = api.util_wavelet(nt, dt, fmax)
    wo, tlo = O.wavelet(nt, dt, fmax)
    assert tl == tlo == tlag
    # independent FFTs in double, both rounded to float: within a few float ulps
    assert np.max(np.abs(w - wo)) <= 4e-7 * np.max(np.abs(wo))


def test_wavelet_peak_frequency_is_fmax_over_3():
    nt, dt, fmax = 4001, 1e-3, 30.0
    r, _ = O.ricker(nt, dt, fmax)
    spec = np.abs(np.fft.rfft(r))
    f = np.fft.rfftfreq(nt, dt)
    assert abs(f[np.argmax(spec)] - fmax / (3 * np.sqrt(np.pi)) * np.sqrt(np.pi)) < 1.0


# ---- damping and indices ----------------------------------------------------------------------
def test_fdm_coefficients_are_the_exact_fractions():
    fdm = [0.001785714285, 0.025396825396, 0.2, 1.6, 2.847222222222]
    exact = [1 / 560, 8 / 315, 1 / 5, 8 / 5, 205 / 72]
    assert max(abs(a - b) for a, b in zip(fdm, exact)) < 1e-11
    # consistency: the Laplacian annihilates constants
    assert abs(2 * (-fdm[0] + fdm[1] - fdm[2] + fdm[3]) - fdm[4]) < 1e-11


@pytest.mark.parametrize("nb,f", [(51, 0.004), (100, 0.004), (21, 0.01)])
def test_b1d_bit_exact(nb, f):
    assert np.array_equal(api.util_b1d(nb, f), O.b1d(nb, f))


def test_grid_indices_bit_exact():
    rng = np.random.default_rng(1)
    c = np.concatenate([rng.uniform(0, 17000, 5000), np.arange(0, 1000, 2.5), [4.99999, 5.0, 5.00001, 14.99]])
    for dh, nb in [(10.0, 100), (25.0, 51), (12.5, 3)]:
        assert np.array_equal(api.util_grid_index(c, dh, nb), O.indices(c, dh, nb))
    # the reference's rounding rule int((c + dh/2)/dh) + nb
    assert list(api.util_grid_index(np.array([0, 4.9, 5.0, 15.0, 24.99]), 10.0, 0)) == [0, 0, 1, 2, 2]


# ---- seeded random-boundary generator -----------------------------------------------------------
def test_ppnd16_matches_scipy():
    p = np.concatenate([np.linspace(1e-6, 1 - 1e-6, 4001), [1e-300, 1e-30, 1e-12, 0.075, 0.925, 1 - 1e-12]])
    ours = np.array([O._lib().orc_ppnd16(float(v)) for v in p])
    ref = ndtri(p)
    assert np.max(np.abs(ours - ref) / np.maximum(1, np.abs(ref))) < 1e-14


def test_det_exp_log():
    x = -np.linspace(0, 700, 3001)
    e = np.array([O._lib().orc_exp(float(v)) for v in x])
    assert np.max(np.abs(e - np.exp(x)) / np.exp(x)) < 1e-15
    y = np.geomspace(1e-300, 1.0, 2001)
    lg = np.array([O._lib().orc_log(float(v)) for v in y])
    assert np.max(np.abs(lg - np.log(y))) < 1e-12


def test_normals_bit_exact_product_vs_oracle():
    for seed in (0, 12345, 2**63 + 11):
        for shot in (0, 3, 80):
            for stream in (1, 2):
                for ctr in list(range(300)) + [10**9, 2**40 + 7]:
                    assert api.util_normal(seed, shot, stream, ctr) == O.normal(seed, shot, stream, ctr)


def test_normals_are_standard_normal():
    v = np.array([O.normal(9, 0, 1, k) for k in range(20000)])
    assert abs(v.mean()) < 0.03 and abs(v.std() - 1) < 0.03


@pytest.mark.parametrize("nzz,nxx,nb,dh,ratio,var,seed,shot", [
    (351, 701, 100, 10.0, 200.0, 500.0, 0, 0), (351, 701, 100, 10.0, 200.0, 500.0, 0, 7),
    (88, 136, 20, 10.0, 60.0, 300.0, 5, 1), (501, 1901, 100, 10.0, 200.0, 1000.0, 42, 3)])
def test_bumps_bit_exact(nzz, nxx, nb, dh, ratio, var, seed, shot):
    a = api.util_bumps(nxx, nzz, nb, dh, ratio, var, seed, shot)
    b = O.bumps(nxx, nzz, nb, dh, ratio, var, seed, shot)
    assert a.shape == b.shape and a.shape[0] > 0
    assert np.array_equal(a, b)
    fnb = nb * dh
    xm, zm = (nxx - 1) * dh, (nzz - 1) * dh
    inner = (a[:, 0] > 0.5 * fnb) & (a[:, 0] < xm - 0.5 * fnb) & (a[:, 1] > 0.5 * fnb) & (a[:, 1] < zm - 0.5 * fnb)
    assert not inner.any()
    assert np.all((a[:, 2] >= 0.2 * ratio) & (a[:, 2] <= ratio))
    assert np.all((a[:, 3] >= 0.5 * var) & (a[:, 3] <= var))
    assert set(np.unique(a[:, 4])) <= {-1.0, 1.0}


def test_poisson_disk_minimum_distance():
    b = O.bumps(351, 701, 100, 10.0, 200.0, 500.0, 3, 0)
    # poissonDiskSampling (admin.cpp:172-199) tests only the 3x3 neighbouring cells of size
    # r/sqrt(2), so points keep at least r/sqrt(2) apart (not r)
    d = np.sqrt(((b[:, None, :2] - b[None, :, :2]) ** 2).sum(-1))
    d[np.arange(len(b)), np.arange(len(b))] = np.inf
    assert d.min() >= 200.0 / np.sqrt(2.0) * (1 - 1e-6)


def test_rbc_oracle_structure():
    """random_boundary_bg + gp: interior untouched except rows/cols nb and n-1-nb, clamp respected."""
    rng = np.random.default_rng(0)
    nz, nx, nb, dh = 30, 50, 10, 10.0
    model = rng.uniform(1500, 3000, (nz, nx)).astype(np.float32)
    base = O.expand(model, nb)
    nzz, nxx = base.shape
    bt = O.bumps(nxx, nzz, nb, dh, 40.0, 400.0, 1, 0)
    out = O.rbc(base, nb, dh, 400.0, float(model.min()), float(model.max()), 1, 0, bt)
    assert np.array_equal(out[nb + 1:-nb - 1, nb + 1:-nb - 1], base[nb + 1:-nb - 1, nb + 1:-nb - 1])
    assert out.max() <= model.max() + 400.0 and out.min() >= model.min() - 400.0
    assert not np.array_equal(out[:nb], base[:nb])
