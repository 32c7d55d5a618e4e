"""The benchmark's reference arm (`bench.py --impl reference`).

It must time the reference's own CPU step (main.cpp:93-108 over cpu.cpp and
Two-phase/two-phase.cpp, built unmodified into oracle/_ref) on the same grid
as the GPU arm, and load nothing of this repository's package or oracle
library into its process.
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

REF = os.path.join(ROOT, "oracle", "_ref", "capaz_ref_2ph")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference CPU binaries not built")

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--grid", "24", "20", "12", "--steps", "2", "--warmup", "1"]
sys.path.insert(0, {root!r})
import bench
bench.main()
loaded = [m for m in sys.modules if m.startswith("capaz_b200") or m.startswith("oracle")]
maps = open("/proc/self/maps").read()
print(json.dumps({{"modules": loaded, "so": [s for s in ("libcapaz_b200", "libcapaz_oracle") if s in maps]}}))
"""


def test_reference_arm_is_clean_and_on_the_workload_grid():
    res = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], capture_output=True, text=True,
                         cwd=ROOT, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(ln) for ln in res.stdout.splitlines() if ln.startswith("{")]
    line, probe = lines[0], lines[1]
    assert probe["modules"] == [] and probe["so"] == [], probe
    assert line["impl"] == "reference" and line["value"] > 0 and line["finite"]
    assert line["steps"] == 2 and line["warmup"] == 1
    sys.path.insert(0, ROOT)
    import bench
    # the same config object the GPU arm prints for this grid
    assert line["config"] == bench.workload_config([24, 20, 12], 1)
    assert line["config"]["grid_ref"] == [24, 12, 20]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_ini_is_read_by_the_reference_as_written():
    """The arm's defines.ini gives the reference the workload's fluids: the
    harness reports the grid it read, and a step from the reference's own
    initial state stays finite."""
    sys.path.insert(0, ROOT)
    import bench
    r = bench.reference_cpu_step((20, 16, 10), 3)
    assert r["cells"] == 20 * 16 * 10 and r["finite"] and r["seconds"] > 0
