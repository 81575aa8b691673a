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


def test_layout_stress_of_a_perfect_layout_is_zero():
    """Stress at the best scale: zero for a path laid out on a line (graph
    distance = Euclidean distance up to scale), positive once it is bent."""
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    V = 50
    a = np.arange(V - 1, dtype=np.uint32)
    b = a + 1
    row, col = bench.csr_numpy(V, a, b)
    line = np.stack([3.0 * np.arange(V), np.zeros(V)], 1).reshape(-1)
    assert abs(bench.layout_stress(row, col, line, sources=5)) < 1e-12
    bent = np.stack([np.cos(np.arange(V) * 0.3), np.sin(np.arange(V) * 0.3)], 1).reshape(-1)
    assert bench.layout_stress(row, col, bent, sources=5) > 1e-3


def test_vector_error_definitions():
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    b = np.array([[1.0, 0.0], [0.0, 2.0]])
    a = np.array([[1.1, 0.0], [0.0, 2.0]])
    e = bench.vector_error(a, b)
    assert abs(e["rms_err"] - 0.1 / np.sqrt(5.0)) < 1e-12
    assert abs(e["max_rel_err_per_vertex"] - 0.1) < 1e-12
    assert abs(e["rms_rel_err_per_vertex"] - np.sqrt(0.01 / 2)) < 1e-12
