"""What the trained CNN preconditioner gains over plain FWI (GPU).

A small version of the experiment of `python -m fwi2d_b200.precond`: pairs
made by the FD engine on seeded dipping-layer models, the U-Net trained on
them with the project's kernels, then FWI of a held-out model from the same
1-D start, plain and CNN-preconditioned (fallback to the gradient when the
line search along the network's direction does not cut the misfit).  The
network must cut the data misfit faster than the gradient does, and it must
reach a lower model error than the plain run reaches, in less wall time (the
quantity the preconditioner is judged on: model RMS error against time).  The
training models are held out from the test model (different seeds)."""
import numpy as np
import pytest

from fwi2d_b200 import api, cnn, precond

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SETUP = precond.PairSetup(nz=96, nx=192, nt=1001, nshots=5, nrec=96, boundary=190.0)


@pytest.fixture(scope="module")
def trained(tmp_path_factory):
    root = tmp_path_factory.mktemp("precond")
    X, T = precond.make_pairs(root / "pairs", models=32, stages=3, setup=SETUP, log=None)
    net = cnn.UNet(seed=0)
    hist = precond.train(net, X, T, SETUP, epochs=20, batch=4, lr=1e-3, val=12, log=None)
    return root, net, hist


def test_training_converges(trained):
    _, _, hist = trained
    assert hist["train"][-1] < 0.75 * hist["train"][1]  # epoch 1 starts from the random init
    assert np.isfinite(hist["val"][-1]) and hist["val"][-1] < hist["val"][0]


def test_cnn_direction_cuts_misfit_faster(trained):
    root, net, _ = trained
    vt = precond.true_model(SETUP, 7)
    vs = precond.start_model(vt, SETUP.dh)
    case = precond.write_setup(root / "test", SETUP, vt)
    runs = {}
    for mode in ("plain", "cnn"):
        with api.Context(case.params, api.MODE_INVERSION) as ctx:
            d = ctx.dims
            seis = torch.empty(d.nsrc * d.nrec * d.nt, dtype=torch.float32, device="cuda")
            ctx.model_survey_dev(seis.data_ptr())  # observed data in the true model
            ctx.set_model(vs)
            ctx.set_observed_dev(seis.data_ptr())
            ctx.set_seed(7)
            runs[mode] = precond.fwi(ctx, vt, 3, net if mode == "cnn" else None, log=None)
    plain, cnn_run = runs["plain"], runs["cnn"]
    assert cnn_run.residuo[0] == plain.residuo[0]  # same start
    assert "cnn" in cnn_run.direction
    # residuo[k] is the misfit before update k + 1: compare after two updates
    assert cnn_run.residuo[-1] < plain.residuo[-1], (cnn_run.residuo, plain.residuo)
    assert all(np.isfinite(cnn_run.model_error))
    # model error against wall time: the CNN run gets below the plain run's
    # best error, and gets there before the plain run has finished
    best_plain = min(plain.model_error)
    t_cnn = precond.time_to_error(cnn_run, best_plain * 0.999)
    print(f"\n[precond] model error plain {plain.model_error} ({plain.seconds[-1]:.2f} s), "
          f"cnn {cnn_run.model_error} ({cnn_run.seconds[-1]:.2f} s)")
    assert t_cnn is not None, (plain.model_error, cnn_run.model_error)
    assert t_cnn < plain.seconds[-1], (t_cnn, plain.seconds)


def test_pairs_along_the_network_trajectory(trained):
    """make_pairs given a network steps each stage along the network's direction
    (with the gradient fallback): finite inputs, targets normalised to max 1."""
    root, net, _ = trained
    X, T = precond.make_pairs(root / "follow", models=2, stages=2, setup=SETUP, log=None, net=net)
    assert X.shape[0] == 4 and T.shape[0] == 4
    assert bool(torch.isfinite(X.float()).all()) and bool(torch.isfinite(T).all())
    for k in range(4):
        assert abs(float(T[k].abs().max()) - 1.0) < 1e-6


def test_training_models_are_held_out():
    """The pairs come from seeds TRAIN_SEED0 .. TRAIN_SEED0 + models - 1; the
    FWI test models (seeds 7 and 11 here, the 301 x 1701 model of seed 2 in
    the survey experiment) are none of them."""
    for seed in (2, 7, 11):
        assert not (precond.TRAIN_SEED0 <= seed < precond.TRAIN_SEED0 + 4096)
