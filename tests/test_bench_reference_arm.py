"""The reference arm of bench.py must not load this library.

`bench.py --impl reference` times the reference's own das; its process may map
oracle/ libraries only.  The workload generators it needs are loaded from
their file (bench.workloads()), so the ffdas_b200 package -- whose import
loads libffdas_b200.so -- is never imported.  Checked in a fresh interpreter.
"""
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import sys
sys.path.insert(0, {root!r})
import bench
W = bench.workloads()
wl = W.plane2d(scale=0.1)
assert wl["x"].shape[-1] > 0
from oracle import reference, oracle  # noqa: F401
bad = sorted(m for m in sys.modules if m == "ffdas_b200" or m.startswith("ffdas_b200."))
assert not bad, bad
with open("/proc/self/maps") as f:
    assert "libffdas_b200.so" not in f.read()
print("ok")
"""


def test_reference_arm_imports_do_not_load_the_library():
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT))], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
