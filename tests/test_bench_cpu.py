"""bench.py pieces that run without a GPU: the reference arm's JSON line (the
CPU restatement of the reference path on a sample of the workload) and the
clock sampler's timed-window filter."""
import datetime
import json
import os
import subprocess
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Runs the reference arm in this interpreter, then prints which shared
# objects of the repository the process mapped.
_RUN_AND_LIST_MAPS = """
import runpy, sys
sys.argv = sys.argv[1:]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
with open("/proc/self/maps") as fh:
    libs = sorted({l.split()[-1] for l in fh if l.rstrip().endswith(".so")})
print("MAPPED " + " ".join(x for x in libs if "nrg" in x.rsplit("/", 1)[-1] or "oracle" in x.rsplit("/", 1)[-1]))
"""


@pytest.mark.parametrize("field", ["flame", "ignition"])
def test_reference_arm_json_line(field):
    r = subprocess.run([sys.executable, "-c", _RUN_AND_LIST_MAPS, "bench.py", "--impl", "reference",
                        "--field", field, "--steps", "1", "--warmup", "0", "--cpu-seconds", "0.2"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.strip().splitlines()
    mapped = out[-1].split()[1:]
    # the reference arm runs the oracle only: no library of the product is mapped
    assert any(m.endswith("oracle/liboracle.so") for m in mapped), mapped
    assert not any("libnrg_chem" in m for m in mapped), mapped
    line = json.loads(out[-2])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "cell-updates/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert ("flame field" if field == "flame" else "ignition field") in line["config"]["workload"]


def test_clock_sampler_keeps_the_timed_window():
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0)
    now = time.time()

    def row(t, mhz, cap):
        ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        return [ts, "0", str(mhz), "1965", "900", "0x0", "Not Active", "Not Active", "Not Active",
                "Active" if cap else "Not Active"]

    c.rows = [row(now - 1.0, 1200, False), row(now + 0.1, 1965, True), row(now + 0.3, 1950, False),
              row(now + 5.0, 345, False), ["garbage"]]
    c.t0, c.t1 = now, now + 1.0
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == pytest.approx(1957.5) and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
