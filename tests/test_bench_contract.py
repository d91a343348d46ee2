"""bench.py's roofline traffic comes from a committed ncu capture, and says so (CPU).

roofline.traffic is the DRAM bytes of one launch of the forward variant the
autotuner chose, read from the `dram_bytes_per_launch[<variant>]` line of a
profiles/ summary.  A variant with no committed capture must be reported as
missing (null with the reason), never silently."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_traffic_of_the_resident_kernel_names_its_capture():
    value, source = bench.traffic_from_profiles("resident W=56 IPT=4 grid=143 | us/step: resident=6.0")
    assert value is not None and value > 0
    assert "profiles/fwd_res_kernel_modeling_survey.md" in source


def test_traffic_of_an_uncaptured_variant_is_reported_missing(capsys):
    value, source = bench.traffic_from_profiles("tma T=2 TX=16 S=2 grid=296 | us/step: tma2,16,2=10.0")
    assert value is None
    assert source.startswith("missing")
    assert "roofline.traffic is null" in capsys.readouterr().err
