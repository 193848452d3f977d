"""CPU test of bench.py's reference arm (`--impl reference`): on the small
20^3 workload it prints one JSON line with the fields of the bench contract,
its per-slice counts and slice ends are the reference build's own run of the
workload (tests/golden/pipelines.json), and the process runs the reference's
own code only -- this library's shared object is never loaded."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT, golden

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libpevsl_ref.so")

WRAPPER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "lap20_5slices",
            "--steps", "1", "--warmup", "3"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED", "libpevsl_b200" in maps, "libpevsl_ref" in maps)
"""


@pytest.mark.slow
def test_reference_arm_contract_and_isolation():
    if not os.path.exists(REF_SO):
        pytest.skip("reference build not available")
    p = subprocess.run([sys.executable, "-c", WRAPPER], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["unit"] == "eigenpairs/s"
    assert out["higher_is_better"] is True and out["steps"] == 1 and out["warmup"] >= 3
    assert out["value"] > 0 and out["cpu_baseline"]["kind"] == "reference"
    assert out["cpu_baseline"]["value"] == out["value"] and out["cpu_baseline"]["cores"] >= 1
    assert out["e2e"] == {"value": out["value"], "unit": "eigenpairs/s",
                          "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert out["config"]["workload"] == "lap20_5slices"
    # the extrapolation uses the reference build's own run of the workload
    g = golden("pipelines.json")["lap20_lantr_gauss"]
    assert out["config"]["slice_ends"] == g["sli"]
    assert out["config"]["filter_degree_per_slice"] == g["deg"]
    assert out["config"]["lanczos_steps_per_slice"] == g["its"]
    assert out["config"]["nev_per_slice"] == g["nev"]
    loaded = [ln for ln in p.stdout.splitlines() if ln.startswith("LOADED")]
    assert loaded == ["LOADED False True"]


def test_reference_arm_fits_the_drivers_step_counts():
    """The reference arm's per-step sample shrinks with the step count so the
    whole arm stays near three minutes of sampling: 20 s per step for the
    default few steps, about 7 s at the driver's 5 + 20, never under 2 s."""
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reference_sample_seconds(3, 1) == 20.0
    assert abs(bench.reference_sample_seconds(5, 20) - 7.2) < 1e-12
    assert bench.reference_sample_seconds(50, 200) == 2.0
    for w, k in ((3, 1), (5, 20), (10, 100)):
        assert (w + k) * bench.reference_sample_seconds(w, k) <= 200.0 + 1e-9 or \
            bench.reference_sample_seconds(w, k) == 2.0
