"""Graph files straight to CSR (gvizCudaLoadEdgesFile / gvizCudaLoadObjFile)
against gviz's own loaders (src/utils/graphLoader.c, the reference compiled
from its sources) followed by its adjacency order: the same vertex numbering,
the same neighbour lists, the same failures."""
import numpy as np
import pytest

EDGES_CASES = {
    "plain_1based": "1 2\n2 3\n3 1\n",
    "zero_based_weights_comments": "% header comment\n0 5 0.5\n5 7 1\n\n  % indented comment\n7 0 2\n",
    "duplicates_selfloops": "4 4\n1 2\n2 1\n1 2\n9 4\n",
    "sparse_ids_crlf": "1000000 3\r\n3 77\r\n77 1000000\r\n4000000 3\r\n",
    "tabs_and_blanks": "\t10\t11\n\n11   12\t9.5\n",
    "header": "3 2\n1 2\n2 3\n",
}
EDGES_BAD = {
    "negative": "1 2\n-3 4\n",
    "one_column": "1 2\n3\n",
    "word": "a b\n",
    "empty": "",
    "only_comments": "% nothing\n%\n",
}
OBJ_CASES = {
    "quad_and_tri": "# mesh\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\nf 1 3 2\n",
    "slashes_negative": "v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\nf 1/1/1 2/1/1 3/1/1\n"
                        "v 1 1 0\nf -1//1 -2//1 -3//1\n",
    "shared_edges_isolated": "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 5 5 5\n"
                             "f 1 2 3\nf 3 2 4\nf 4 3 1\ng group\nusemtl m\ns off\n",
    "degenerate": "v 0 0 0\nv 1 0 0\nf 1 1 2\nf 2\nf 1 2\n",
}
OBJ_BAD = {"zero_index": "v 0 0 0\nf 0 1\n", "out_of_range": "v 0 0 0\nf 1 2\n",
           "no_vertices": "# empty\n", "bad_token": "v 0 0 0\nv 1 1 1\nf 1 x\n"}


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return p


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("case", sorted(EDGES_CASES))
def test_edges_file_matches_gviz(ref, tmp_path, case, directed):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".edges", EDGES_CASES[case])
    skip = case == "header"
    want = ref.load_edges_csr(p, directed, skip)
    row, col, ext = graphs.load_edges_file(p, directed, skip)
    assert want is not None
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])
    assert len(ext) == len(row) - 1


def test_edges_file_external_ids(ref, tmp_path):
    """Ids far apart: gviz's loader sizes its id map by max - min + 1 and
    cannot allocate it here; this loader maps only the ids present."""
    from grapher_b200 import graphs
    p = _write(tmp_path, "ids.edges", "1000000 3\n3 77\n77 1000000\n5000000000 3\n")
    row, col, ext = graphs.load_edges_file(p)
    assert ext.tolist() == [1000000, 3, 77, 5000000000]
    assert row.tolist() == [0, 2, 5, 7, 8]
    assert col.tolist() == [1, 2, 0, 2, 3, 1, 0, 1]


@pytest.mark.parametrize("case", sorted(EDGES_BAD))
def test_edges_file_failures_match_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".edges", EDGES_BAD[case])
    assert ref.load_edges_csr(p) is None
    with pytest.raises(OSError):
        graphs.load_edges_file(p)


def test_missing_file(tmp_path):
    from grapher_b200 import graphs
    with pytest.raises(OSError):
        graphs.load_edges_file(tmp_path / "absent.edges")
    with pytest.raises(OSError):
        graphs.load_obj_file(tmp_path / "absent.obj")


@pytest.mark.parametrize("case", sorted(OBJ_CASES))
def test_obj_file_matches_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".obj", OBJ_CASES[case])
    want = ref.load_obj_csr(p)
    row, col = graphs.load_obj_file(p)
    assert want is not None
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])


@pytest.mark.parametrize("case", sorted(OBJ_BAD))
def test_obj_file_failures_match_gviz(ref, tmp_path, case):
    from grapher_b200 import graphs
    p = _write(tmp_path, case + ".obj", OBJ_BAD[case])
    assert ref.load_obj_csr(p) is None
    with pytest.raises(OSError):
        graphs.load_obj_file(p)


def test_random_edges_file_matches_gviz(ref, tmp_path):
    """A seeded 200k-line file with duplicates, self-loops and scattered ids."""
    from grapher_b200 import graphs
    rng = np.random.default_rng(5)
    ids = rng.choice(10 ** 7, 30000, replace=False) + 1
    u = ids[rng.integers(0, len(ids), 200000)]
    v = ids[rng.integers(0, len(ids), 200000)]
    lines = "\n".join(f"{a} {b}" for a, b in zip(u, v))
    p = _write(tmp_path, "rand.edges", "% random\n" + lines + "\n")
    want = ref.load_edges_csr(p)
    row, col, ext = graphs.load_edges_file(p)
    assert np.array_equal(row, want[0]) and np.array_equal(col, want[1])
    assert ext[0] == u[0]
