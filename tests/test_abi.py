"""The C-ABI library loads and exports every function the headers in include/ declare."""
import ctypes
import re
from pathlib import Path

from fwi2d_b200 import api

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))


def declared_functions() -> set[str]:
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(fwi_\w+)\s*\(", text))
    return names


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("fwi_ctx_create", "fwi_model_shot", "fwi_rtm_shot", "fwi_compute_gradient", "fwi_linesearch_trial",
                 "fwi_update_model", "fwi_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(api.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    assert declared_functions() == set(api.SIGNATURES)


def test_executables_built():
    from fwi2d_b200 import build as b
    for app in b.APPS:
        assert (b.BIN / app).exists()


def test_create_failure_reports_error_without_gpu(tmp_path):
    # a missing parameters file fails before any CUDA call
    try:
        api.Context(tmp_path / "nope.txt", api.MODE_MODELING)
    except api.FwiError as e:
        assert e.code == -2 and "could not be opened" in str(e)
    else:
        raise AssertionError("expected FwiError")


def test_nn_kernels_refuse_unsupported_sizes_without_gpu():
    """The CNN entry points check sizes and alignment before any CUDA call:
    channel counts that are not multiples of 8 (16 for the convolutions),
    buffers off a 16-byte boundary and ReLU-gradient lengths that are not
    multiples of 8 return FWI_ERR_ARG (-8)."""
    L = api.lib()
    ok, odd = 1 << 20, (1 << 20) + 8  # addresses only compared, never read
    assert L.fwi_nn_pool2(ok, 1, 4, 4, 12, ok, None) == -8
    assert L.fwi_nn_pool2(odd, 1, 4, 4, 16, ok, None) == -8
    assert L.fwi_nn_pool2_bwd(ok, 1, 4, 4, 20, ok, 0, None) == -8
    assert L.fwi_nn_upcat(ok, 2, 2, 12, ok, 1, 4, 4, 16, ok, None) == -8
    assert L.fwi_nn_upcat(ok, 2, 2, 16, ok, 1, 4, 4, 16, odd, None) == -8
    assert L.fwi_nn_upcat_bwd(ok, 1, 4, 4, 16, 4, 2, 2, ok, 0, ok, 0, None) == -8
    assert L.fwi_nn_relu_bwd(ok, ok, 100, ok, None) == -8
    assert L.fwi_nn_relu_bwd(ok, odd, 128, ok, None) == -8
    assert L.fwi_nn_mse(ok, 12, ok, None, 16, 1.0, ok, ok, ok, None) == -8
    assert L.fwi_nn_conv3x3(ok, 1, 8, 8, 24, ok, None, 16, 0, ok, None, None) == -8
    assert L.fwi_nn_conv3x3(odd, 1, 8, 8, 16, ok, None, 16, 0, ok, None, None) == -8
    assert L.fwi_nn_conv3x3(ok, 1, 8, 8, 16, ok, None, 272, 0, ok, None, None) == -8
