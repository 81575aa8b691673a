"""CPU checks of libgvizcuda: it loads, exports every entry point its headers
declare, and its host helpers reproduce the reference's fixture graphs and
initial placement (no kernel runs here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gvizCuda\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from grapher_b200 import _native
    lib = _native.lib()
    names = _declared("gvizcuda.h")
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_workloads_library_exports_its_header_and_stays_apart():
    """libgvizworkloads exports include/gvizworkloads.h, and it does not pull
    in libgvizcuda (the CPU reference timing builds its graphs with it)."""
    import subprocess
    from grapher_b200 import _native
    lib = _native.workloads_lib()
    names = [n for n in re.findall(r"\b(gvizGen\w+)\s*\(",
                                   re.sub(r"/\*.*?\*/", "",
                                          open(os.path.join(ROOT, "include",
                                                            "gvizworkloads.h")).read(),
                                          flags=re.S))]
    assert len(names) == 5
    assert all(hasattr(lib, n) for n in names)
    assert set(names) <= set(_native._WSIGS)
    deps = subprocess.run(["ldd", _native.WORKLOADS_PATH], capture_output=True,
                          text=True).stdout
    assert "gvizcuda" not in deps and "libcuda" not in deps and "cudart" not in deps


def test_glue_library_exports_its_headers():
    """The gviz-side glue (built only where gviz's headers are) exports every
    entry point of include/gvizCudaForceEmbedder.h and gvizCudaGripEmbedder.h."""
    import subprocess
    glue = os.path.join(ROOT, "grapher_b200", "lib", "libgvizcuda_gviz.so")
    if not os.path.exists(glue):
        pytest.skip("gviz glue not built here")
    out = subprocess.run(["nm", "-D", "--defined-only", glue], capture_output=True,
                         text=True).stdout
    defined = set(line.split()[-1] for line in out.splitlines() if line.strip())
    for header in ("gvizCudaForceEmbedder.h", "gvizCudaGripEmbedder.h"):
        missing = [n for n in _declared(header) if n not in defined]
        assert not missing, (header, missing)


def test_python_binding_covers_the_header():
    from grapher_b200 import _native
    names = set(_declared("gvizcuda.h"))
    assert names <= set(_native._SIGS), sorted(names - set(_native._SIGS))


def test_grid_matches_reference_fixture():
    from grapher_b200 import graphs
    g = golden("traj_grid32_fr_theta05")
    a, b = graphs.grid(32, 32)
    assert np.array_equal(a, g["ea"]) and np.array_equal(b, g["eb"])


@pytest.mark.parametrize("name,args", [("traj_rc300_linlog_theta08_grav_overlap", (300, 0.02, 5)),
                                       ("traj_rc200_fr_exact", (200, 0.05, 9)),
                                       ("traj_rc500_linlog_theta12_k3", (500, 0.0, 3))])
def test_random_connected_matches_reference_fixture(name, args):
    from grapher_b200 import graphs
    g = golden(name)
    a, b = graphs.random_connected(*args)
    assert np.array_equal(a, g["ea"]) and np.array_equal(b, g["eb"])


def test_randomize_positions_matches_reference_begin():
    # Begin(seed) draws x then y per vertex with rand_r
    # (src/embedders/gvizEmbeddedGraph.c:406-426)
    from grapher_b200 import graphs
    g = golden("traj_grid32_fr_theta05")
    xy = graphs.randomize_positions(1024, 1.0, int(g["seed"]))
    assert np.array_equal(xy, g["x0"])


def test_csr_follows_add_edge_order():
    from grapher_b200 import graphs
    row, col = graphs.to_csr(4, np.array([0, 2, 1, 3], np.uint32), np.array([1, 0, 1, 0], np.uint32))
    # (1,1) is a self loop: appended twice to vertex 1's list
    assert row.tolist() == [0, 3, 6, 7, 8]
    assert col.tolist() == [1, 2, 3, 0, 1, 1, 0, 0]


def test_barabasi_albert_shape():
    from grapher_b200 import graphs
    a, b = graphs.barabasi_albert(5000, 4, 7)
    assert len(a) == 4 * 5000 - 10
    assert np.all(a != b)
    keys = np.minimum(a, b).astype(np.uint64) << 32 | np.maximum(a, b)
    assert len(np.unique(keys)) == len(keys)
    deg = np.bincount(np.concatenate([a, b]), minlength=5000)
    assert deg.min() >= 4 and deg.max() > 100  # preferential attachment hubs


def test_erdos_renyi_and_rmat():
    from grapher_b200 import graphs
    a, b = graphs.erdos_renyi(1000, 4000, 3)
    assert len(a) == 4000 and np.all(a != b)
    keys = np.minimum(a, b).astype(np.uint64) << 32 | np.maximum(a, b)
    assert len(np.unique(keys)) == 4000
    a, b = graphs.rmat(10, 8000, seed=5)
    assert np.all(a < b) and len(a) < 8000
    keys = a.astype(np.uint64) << 32 | b
    assert len(np.unique(keys)) == len(keys)


def test_generators_are_deterministic():
    from grapher_b200 import graphs
    for f, args in [(graphs.barabasi_albert, (3000, 4, 1)), (graphs.erdos_renyi, (500, 900, 2)),
                    (graphs.rmat, (9, 2000, 0.57, 0.19, 0.19, 4))]:
        a1, b1 = f(*args)
        a2, b2 = f(*args)
        assert np.array_equal(a1, a2) and np.array_equal(b1, b2)


def test_create_without_device_fails_loudly():
    from grapher_b200 import ForceLayout, GvizCudaError, graphs
    from grapher_b200 import _native
    n = ctypes.c_int()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    a, b = graphs.grid(3, 3)
    row, col = graphs.to_csr(9, a, b)
    with pytest.raises(GvizCudaError) as e:
        ForceLayout(row, col)
    assert e.value.code == -8  # GVIZ_CUDA_ERR_NO_DEVICE
    assert _native.lib().gvizCudaErrorString(-8) == b"no usable CUDA device"
    del n
