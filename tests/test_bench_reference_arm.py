"""The benchmark's reference arm (`bench.py --impl reference`) on the host:
the reference's own build_tree (oracle/_ref/ref_driver, compiled from the
reference sources) times a small RMAT build and prints one JSON line with the
contract's keys, without importing this package (its input is generated by
the driver itself), so the reference arm's number owes nothing to the
product library.  CPU only."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

PROBE = """
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--scale", "12", "--steps", "2", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
print(json.dumps({"package_imported": any(m == "risgraph_b200" or m.startswith("risgraph_b200.")
                                          for m in sys.modules)}))
"""


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference-built oracle is not built here")
def test_reference_arm_prints_the_contract_line_without_the_package():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 2, out.stdout
    line, probe = lines
    assert probe["package_imported"] is False
    assert line["impl"] == "reference" and line["unit"] == "GTEPS" and line["value"] > 0
    for k in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "dtype",
              "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["scale"] == 12
