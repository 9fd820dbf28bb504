"""The bench line's roofline is read from the committed ncu summaries under
profiles/: every benchmark workload has one, its key lines parse, and they
carry the instruction count the issue roof needs (per timed launch, or per
path for the multi-launch wavefront engine). With the timed launch's figures
the roofline object is the issue bound with a fraction below the roof."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

PEAKS = {"hbm_gbs": 6540.5}


@pytest.mark.parametrize("workload", sorted(bench.PROFILE))
def test_profile_keys(workload):
    f = ROOT / "profiles" / bench.PROFILE[workload]
    assert f.exists(), f
    prof = bench.profiled_figures(bench.PROFILE[workload])
    assert prof.get("kernel") and prof.get("ncu_case")
    assert prof.get("inst_executed_per_launch") or prof.get("inst_executed_per_path")
    assert 0.9 <= float(prof.get("kernel_share_of_step", 1.0)) <= 1.0
    # only the key block is read: no prose line parses as a key
    for k in prof:
        assert " " not in k, k


# (workload, timed step ms, live kernel ms, segments, paths, pixels): the
# figures of the bench lines the summaries were captured beside
CASES = [("cornell", 14.88, 14.87, 1.68e8, 67108864, 262144),
         ("one_weekend", 0.80, 0.78, 5.74e6, 2880000, 90000),
         ("icospheres", 27.6, 27.6, 1.97e8, 132710400, 2073600),
         ("sdf_field", 2657.0, None, 3.8e9, 1887436800, 14745600)]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_roofline_is_the_issue_bound(case):
    workload, t_ms, k_ms, segs, paths, npx = case
    r = bench.roofline(workload, PEAKS, "measured", 1965.0, t_ms, k_ms, segs, paths, npx)
    assert r["bound"] == "issue"
    assert 0.3 < r["frac"] < 1.05, r["frac"]
    assert r["peak"] == pytest.approx(148 * 4 * 1.965, rel=1e-6)
