"""The bench's reference arm on the CPU: it prints the same metric string as
the repo's own arm for the same workload, and the process never maps
libgvizcuda (its graphs come from libgvizworkloads, the reference from
oracle/_ref)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'grid32', '--steps', '2',
            '--warmup', '0']
try:
    runpy.run_path('bench.py', run_name='__main__')
except SystemExit:
    pass
maps = open('/proc/self/maps').read()
print('MAPPED', int('libgvizcuda.so' in maps), int('libgviz_ref.so' in maps))
"""


def test_reference_arm_matches_metric_and_leaves_the_library_unloaded():
    sys.path.insert(0, ROOT)
    import bench
    from oracle.bindings import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref not built here")
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    line = json.loads(next(ln for ln in lines if ln.startswith("{")))
    assert line["impl"] == "reference"
    assert line["metric"] == bench.Workload("grid32").metric()
    assert line["cpu_baseline"]["cpu_model"]
    mapped = next(ln for ln in lines if ln.startswith("MAPPED")).split()
    assert mapped[1] == "0", "the reference arm loaded libgvizcuda"
    assert mapped[2] == "1"


def test_learned_metric_is_the_headline_string():
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "BASELINE.json")) as f:
        metric = json.load(f)["metric"]
    w = bench.Workload.__new__(bench.Workload)
    w.name = "ba1m_learned"
    assert w.metric() == metric
