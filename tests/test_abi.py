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
