"""bench.py's reference arm on the CPU: the JSON line the driver reads, and that the arm runs the
oracle without loading this package or any of its native libraries (so its timing is the CPU
reference alone)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    if e.code not in (0, None):
        raise
pkg = sorted(m for m in sys.modules if m == "diff_envshade_b200" or m.startswith("diff_envshade_b200."))
maps = open("/proc/self/maps").read()
native = sorted({l.split()[-1] for l in maps.splitlines() if "libdes_b200" in l or "diff_envshade_b200/_C" in l})
print("CHILD-REPORT", repr(pkg), repr(native))
"""


def test_reference_arm_line_and_isolation():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", _CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    report = [l for l in lines if l.startswith("CHILD-REPORT")]
    assert report, r.stdout[-2000:]
    pkg, native = report[0].split(" ", 2)[1:]
    assert pkg == "[]", f"the reference arm imported the package: {pkg}"
    assert native == "[]", f"the reference arm mapped native code of the package: {native}"
    data = [json.loads(l) for l in lines if l.startswith("{")]
    assert len(data) == 1
    d = data[0]
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["config"]["workload"].startswith("vis-70k")
